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
//   5. group    segmented sums of price per fk over the joined prefix; every
//               row writes a group record, ORCompact moves the groups to the
//               front (public bound: the dimension size)
//   6. top-k    groups ordered on (sum desc, fk asc): for k <= 16 every
//               4096-row tile is sorted in one in-tile pass, its best 16
//               rows are gathered and only those candidates are fully
//               sorted; otherwise a full bitonic sort; first k
// Record layout of the union (2 u64 words):
//   w0 = [63:32] key ^ 0x80000000 | [31] tag (0 dim, 1 fact) | [30] row passes
//        its side's filter | [29] joined (set by fill) ; w1 = price (fact rows)
#include "net_impl.cuh"
#include "segagg.cuh"

namespace velo {

// ties (fact rows of one key) are aggregated, their order is irrelevant; the
// union sorts on the whole of w0, whose bits below the (key, tag) pair only
// refine that order
using JRec = RowRec<2, 1, false, KEY_FULL>;
using GRec = RowRec<3, 1, false>;
using TRec = RowRec<3, 3, false>;
constexpr uint64_t J_KEYTAG = 0xFFFFFFFF80000000ull;
constexpr uint64_t J_JOINED = 1ull << 29;
constexpr int J_LT = 12; // 4096-row tiles (CTA shape per record width: Tile12)
// up to 8 fused global levels: 16 contiguous rows of 8-byte words fill a line
constexpr int J_LMAX = J_LT - 4 < 8 ? J_LT - 4 : 8;
constexpr int J_TOPK_CAND = 16; // candidates kept per sorted tile (k <= 16 takes the tile path)

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

__global__ void __launch_bounds__(FILL_THREADS) k_fill_summary(const uint64_t* w0, DimCarry* tile_last)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_summary"));
    // the tile's last dimension row: every thread keeps the last one of its
    // stride (rows are visited in increasing order), then a max-index
    // reduction picks the overall last
    __shared__ DimCarry sm[FILL_THREADS];
    __shared__ int idx[FILL_THREADS];
    const size_t base = (size_t)blockIdx.x * FILL_TS;
    DimCarry c { 0, 0, 0 };
    int last = -1;
    for (int i = threadIdx.x; i < FILL_TS; i += FILL_THREADS) {
        VELO_TRACE_AT(TS_FILL, w0 + base + i);
        const DimCarry d = dim_of(w0[base + i]);
        c = dim_combine(c, d);
        last = d.has ? i : last;
    }
    sm[threadIdx.x] = c;
    idx[threadIdx.x] = last;
    __syncthreads();
    for (int off = FILL_THREADS / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            const int x = idx[threadIdx.x], y = idx[threadIdx.x + off];
            const bool take_y = y > x;
            sm[threadIdx.x] = take_y ? sm[threadIdx.x + off] : sm[threadIdx.x];
            idx[threadIdx.x] = take_y ? y : x;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        tile_last[blockIdx.x] = sm[0];
}

// exclusive "last dimension row" scan over tiles; one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_fill_carries(const DimCarry* tile_last, int ntiles, DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_carries"));
    __shared__ DimCarry sm[1024];
    const int per = (ntiles + 1023) / 1024;
    const int t0 = threadIdx.x * per, t1 = min(ntiles, t0 + per);
    DimCarry c { 0, 0, 0 };
    for (int t = t0; t < t1; t++) {
        VELO_TRACE_AT(TS_FILL, tile_last + t);
        c = dim_combine(c, tile_last[t]);
    }
    sm[threadIdx.x] = c;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        DimCarry prev = (int)threadIdx.x >= off ? sm[threadIdx.x - off] : DimCarry { 0, 0, 0 };
        __syncthreads();
        sm[threadIdx.x] = dim_combine(prev, sm[threadIdx.x]);
        __syncthreads();
    }
    DimCarry run = threadIdx.x > 0 ? sm[threadIdx.x - 1] : DimCarry { 0, 0, 0 };
    for (int t = t0; t < t1; t++) {
        carry[t] = run;
        run = dim_combine(run, tile_last[t]);
    }
}

__global__ void __launch_bounds__(FILL_THREADS) k_fill_apply(uint64_t* w0, const DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_apply"));
    __shared__ uint64_t sw[FILL_TS];
    __shared__ DimCarry st[FILL_THREADS];
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
    st[threadIdx.x] = mine;
    __syncthreads();
    for (int off = 1; off < FILL_THREADS; off <<= 1) {
        DimCarry prev = (int)threadIdx.x >= off ? st[threadIdx.x - off] : DimCarry { 0, 0, 0 };
        __syncthreads();
        st[threadIdx.x] = dim_combine(prev, st[threadIdx.x]);
        __syncthreads();
    }
    DimCarry run = dim_combine(carry[blockIdx.x], threadIdx.x > 0 ? st[threadIdx.x - 1] : DimCarry { 0, 0, 0 });
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

// ---- group records -> top-k sort records ------------------------------------
// g0 = [63] not a group | [31:0] fk ^ sign ; g1 = sum price ; g2 = count
// t0 = [63] not a group ; t1 = ~(sum ^ sign) (sum descending) ; t2 = fk << 32 | count
__global__ void k_topk_pack(const uint64_t* g0, const uint64_t* g1, const uint64_t* g2, size_t n, uint64_t* t0,
                            uint64_t* t1, uint64_t* t2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_pack"));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, n); i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t a = g0[i];
        t0[i] = a & (1ull << 63);
        t1[i] = ~(g1[i] ^ 0x8000000000000000ull);
        t2[i] = ((a & 0xFFFFFFFFull) << 32) | (g2[i] & 0xFFFFFFFFull);
    }
}

// the best `c` rows of every sorted tile of 2^lt rows: tiles with bit lt of
// their first row clear were sorted ascending (best first), the others
// descending (best last); row positions depend only on the tile index
__global__ void k_topk_candidates(const uint64_t* t0, const uint64_t* t1, const uint64_t* t2, int lt, int c,
                                  size_t ntiles, uint64_t* c0, uint64_t* c1, uint64_t* c2)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_candidates"));
    const size_t total = ntiles * (size_t)c;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; VELO_GRID_COND(i, total);
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t tile = i / (size_t)c, r = i % (size_t)c;
        const size_t base = tile << lt;
        const size_t src = (tile & 1) ? base + ((size_t)1 << lt) - 1 - r : base + r;
        c0[i] = t0[src];
        c1[i] = t1[src];
        c2[i] = t2[src];
    }
}

__global__ void k_topk_out(const uint64_t* t0, const uint64_t* t1, const uint64_t* t2, size_t k, int64_t* out,
                           const uint64_t* n_groups, const uint64_t* n_joined, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_out"));
    for (size_t i = threadIdx.x; i < k; i += blockDim.x) {
        VELO_TRACE_AT(TS_TOPK, t0 + i);
        const bool ok = (t0[i] >> 63) == 0;
        out[i * 3 + 0] = ok ? (int64_t)(int32_t)((uint32_t)(t2[i] >> 32) ^ 0x80000000u) : 0;
        out[i * 3 + 1] = ok ? (int64_t)(~t1[i] ^ 0x8000000000000000ull) : 0;
        out[i * 3 + 2] = ok ? (int64_t)(t2[i] & 0xFFFFFFFFull) : 0;
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

__global__ void __launch_bounds__(SEG_THREADS) k_jseg_emit_rows(JRec::Cols c, int ntiles, const SegTileAgg* aggs,
                                                                const int64_t* carry_in, GRec::Cols g)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_jseg_emit_rows"));
    extern __shared__ __align__(16) char sm[];
    JSeg::emit_rows(c.w, blockIdx.x, ntiles, aggs, carry_in, g.w, JoinAgg::Params {}, sm);
}

struct JoinScratch {
    uint64_t* u[2];      // union records
    uint64_t* g[3];      // group records
    uint64_t* t[3];      // top-k sort records (aliases the union area)
    uint32_t* counts;
    uint32_t* prefix;
    uint64_t* n_joined;
    uint32_t* gcounts;
    uint32_t* gprefix;
    uint64_t* n_grp_rows;
    DimCarry* tile_last;
    DimCarry* fcarry;
    SegTileAgg* aggs;
    int64_t* runs;
    int64_t* carry;
    uint32_t* tail_prefix;
    uint64_t* n_groups;
    size_t bytes, n_rec, n_top;
};

static JoinScratch join_layout(char* base, size_t nd, size_t nf)
{
    JoinScratch s {};
    size_t n_rec = next_pow2(nd + nf);
    const size_t floor_rows = (size_t)1 << J_LT;
    n_rec = n_rec < floor_rows ? floor_rows : n_rec;
    n_rec = n_rec < (size_t)SEG_TS ? (size_t)SEG_TS : n_rec;
    s.n_rec = n_rec;
    s.n_top = next_pow2(nd);
    const size_t ntc = n_rec >> J_LT, nts = n_rec / SEG_TS, ntf = n_rec / FILL_TS;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes, 256);
        return p;
    };
    for (int i = 0; i < 2; i++)
        s.u[i] = reinterpret_cast<uint64_t*>(take(n_rec * 8));
    for (int i = 0; i < 3; i++)
        s.g[i] = reinterpret_cast<uint64_t*>(take(n_rec * 8));
    s.counts = reinterpret_cast<uint32_t*>(take(ntc * 4));
    s.prefix = reinterpret_cast<uint32_t*>(take((ntc + 1) * 4));
    s.n_joined = reinterpret_cast<uint64_t*>(take(8));
    s.gcounts = reinterpret_cast<uint32_t*>(take(ntc * 4));
    s.gprefix = reinterpret_cast<uint32_t*>(take((ntc + 1) * 4));
    s.n_grp_rows = reinterpret_cast<uint64_t*>(take(8));
    s.tile_last = reinterpret_cast<DimCarry*>(take(ntf * sizeof(DimCarry)));
    s.fcarry = reinterpret_cast<DimCarry*>(take(ntf * sizeof(DimCarry)));
    s.aggs = reinterpret_cast<SegTileAgg*>(take(nts * sizeof(SegTileAgg)));
    s.runs = reinterpret_cast<int64_t*>(take(nts * JoinAgg::V * 8));
    s.carry = reinterpret_cast<int64_t*>(take(nts * JoinAgg::V * 8));
    s.tail_prefix = reinterpret_cast<uint32_t*>(take(nts * 4));
    s.n_groups = reinterpret_cast<uint64_t*>(take(8));
    s.bytes = off;
    // the top-k records reuse the union area (free after the group-by) plus
    // the group area's third word
    s.t[0] = s.u[0];
    s.t[1] = s.u[1];
    s.t[2] = base ? reinterpret_cast<uint64_t*>(base) + 0 : nullptr;
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
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_jseg_emit_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JSeg::SMEM),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_join_groupby_topk_scratch_bytes(size_t n_dim, size_t n_fact)
{
    JoinScratch s = join_layout(nullptr, n_dim, n_fact);
    // the top-k records need a third word array of next_pow2(n_dim) rows
    return s.bytes + align_up(s.n_top * 8, 256);
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
    const size_t need = s.bytes + align_up(s.n_top * 8, 256);
    if (!d_scratch || scratch_bytes < need) {
        set_error("velo_join_groupby_topk: scratch must hold velo_join_groupby_topk_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    s.t[2] = reinterpret_cast<uint64_t*>(static_cast<char*>(d_scratch) + s.bytes);
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
    if (logU > 0) {
        std::vector<NetPass> passes;
        plan_sort(logU, J_LT, J_LMAX, passes);
        rc = launch_net12<JRec>(uc, NetGeom { (size_t)1 << logU, logU, 0 }, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
    }
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
    // compaction keeps the sorted order of the joined rows)
    const int nts = (int)(s.n_rec / SEG_TS);
    GRec::Cols gc;
    for (int i = 0; i < 3; i++) {
        gc.w[i] = s.g[i];
        gc.pad[i] = ~0ull;
    }
    gc.mask[0] = ~0ull;
    gc.mark_bit = 63;
    gc.mark_inv = 1;
    gc.mark_word = 0;
    k_jseg_summary<<<nts, SEG_THREADS, JSeg::SMEM_IN, st>>>(uc, s.aggs, s.runs);
    k_jseg_carries<<<1, 1024, JoinAgg::V * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, nts, s.carry,
                                                                            s.tail_prefix, s.n_groups);
    k_jseg_emit_rows<<<nts, SEG_THREADS, JSeg::SMEM, st>>>(uc, nts, s.aggs, s.carry, gc);
    VELO_CUDA_TRY(cudaGetLastError(), "join group-by launch");
    {
        const int ntc = logR > J_LT ? 1 << (logR - J_LT) : 1;
        k_count_marks<GRec><<<ntc, 256, 0, st>>>(gc, s.n_rec, J_LT, s.gcounts);
        k_scan_tiles<<<1, 1024, 0, st>>>(s.gcounts, ntc, s.gprefix, s.n_grp_rows);
        std::vector<NetPass> passes;
        plan_compact(logR, J_LT, J_LMAX, passes);
        rc = launch_net12<GRec>(gc, NetGeom { s.n_rec, logR, 0 }, passes, s.gprefix, st);
        if (rc != VELO_OK)
            return rc;
    }
    tm.mark();
    // 6. top-k: sort the first next_pow2(n_dim) group records (the public
    // bound on the number of groups) on (sum desc, fk asc)
    const size_t n_top = s.n_top;
    k_topk_pack<<<148 * 4, 256, 0, st>>>(s.g[0], s.g[1], s.g[2], n_top, s.t[0], s.t[1], s.t[2]);
    TRec::Cols tc;
    for (int i = 0; i < 3; i++) {
        tc.w[i] = s.t[i];
        tc.pad[i] = ~0ull;
    }
    tc.mask[0] = 1ull << 63;
    tc.mask[1] = ~0ull;
    tc.mask[2] = 0xFFFFFFFF00000000ull;
    tc.mark_bit = 63;
    tc.mark_inv = 1;
    tc.mark_word = 0;
    const int logT = ilog2_floor(n_top);
    const uint64_t* w0 = s.t[0];
    const uint64_t* w1 = s.t[1];
    const uint64_t* w2 = s.t[2];
    if (logT > J_LT && k <= J_TOPK_CAND) {
        // top-k without a full sort: the in-tile pass sorts every tile of
        // 2^J_LT rows, the best J_TOPK_CAND rows of each tile are gathered
        // (the overall best k lie among them), and the candidates are sorted
        std::vector<NetPass> passes { NetPass { P_SORT_TILE, J_LT, 0, 0 } };
        rc = launch_net12<TRec>(tc, NetGeom { n_top, logT, 0 }, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
        const size_t ntiles = n_top >> J_LT;
        const size_t nc = ntiles * J_TOPK_CAND;
        k_topk_candidates<<<148 * 4, 256, 0, st>>>(s.t[0], s.t[1], s.t[2], J_LT, J_TOPK_CAND, ntiles, s.g[0],
                                                    s.g[1], s.g[2]);
        VELO_CUDA_TRY(cudaGetLastError(), "top-k candidates launch");
        TRec::Cols cc = tc;
        for (int i = 0; i < 3; i++)
            cc.w[i] = s.g[i];
        const int logC = ilog2_floor(nc);
        passes.clear();
        plan_sort(logC, J_LT, J_LMAX, passes);
        rc = launch_net12<TRec>(cc, NetGeom { nc, logC, 0 }, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
        w0 = s.g[0];
        w1 = s.g[1];
        w2 = s.g[2];
    } else if (logT > 0) {
        std::vector<NetPass> passes;
        plan_sort(logT, J_LT, J_LMAX, passes);
        rc = launch_net12<TRec>(tc, NetGeom { n_top, logT, 0 }, passes, nullptr, st);
        if (rc != VELO_OK)
            return rc;
    }
    const size_t kk = k < n_top ? k : n_top;
    k_topk_out<<<1, 256, 0, st>>>(w0, w1, w2, kk, d_out, s.n_groups, s.n_joined, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "top-k launch");
    if (kk < k)
        VELO_CUDA_TRY(cudaMemsetAsync(d_out + kk * 3, 0, (k - kk) * 3 * 8, st), "cudaMemsetAsync");
    tm.mark();
    tm.finish();
    return VELO_OK;
}
