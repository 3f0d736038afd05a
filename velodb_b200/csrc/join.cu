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
#include "join.cuh"

namespace velo {

__global__ void __launch_bounds__(256) k_join_pack(const int32_t* dk, const int32_t* dd, size_t nd, const int32_t* ff,
                                                   const int64_t* fp, size_t nf, int32_t date_hi, int64_t price_hi,
                                                   size_t n_rec, uint64_t* w0, uint64_t* w1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_join_pack"));
    join_pack_body(dk, dd, nd, ff, fp, nf, date_hi, price_hi, n_rec, w0, w1, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(FILL_THREADS) k_fill_summary(const uint64_t* w0, DimCarry* tile_last)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_summary"));
    __shared__ DimCarry sm[FILL_THREADS / 32];
    __shared__ int idx[FILL_THREADS / 32];
    fill_summary_tile(w0, tile_last, blockIdx.x, sm, idx);
}

__global__ void __launch_bounds__(1024) k_fill_carries(const DimCarry* tile_last, int ntiles, DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_carries"));
    __shared__ DimCarry wsm[33];
    fill_carries_body(tile_last, ntiles, carry, wsm);
}

__global__ void __launch_bounds__(FILL_THREADS) k_fill_apply(uint64_t* w0, const DimCarry* carry)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_fill_apply"));
    __shared__ uint64_t sw[FILL_TS_PAD];
    __shared__ DimCarry wsm[33];
    fill_apply_tile(w0, carry, blockIdx.x, sw, wsm);
}

__global__ void __launch_bounds__(TK_RED_THREADS) k_topk_reduce(const uint64_t* in0, const uint64_t* in1, int rn,
                                                                int c, uint64_t* out0, uint64_t* out1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_reduce"));
    extern __shared__ __align__(16) char sm[];
    topk_reduce_tile<TK_RED_ROWS / 2 / TK_RED_THREADS>(in0, in1, rn, c, out0, out1, blockIdx.x, sm);
}

__global__ void k_topk_out(const uint64_t* t0, const uint64_t* t1, size_t k, int64_t* out, const uint64_t* n_groups,
                           const uint64_t* n_joined, uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_topk_out"));
    topk_out_body(t0, t1, k, out, n_groups, n_joined, d_counts);
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

__global__ void __launch_bounds__(SEG_THREADS, 5) k_jseg_emit_topk(JRec::Cols c, int ntiles, const SegTileAgg* aggs,
                                                                const int64_t* carry_in, int cand, uint64_t* out0,
                                                                uint64_t* out1)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_jseg_emit_topk"));
    extern __shared__ __align__(16) char sm[];
    jseg_emit_topk_tile(c, ntiles, aggs, carry_in, cand, out0, out1, blockIdx.x, sm);
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
    const size_t topk_smem = cand == 16 ? JSEG_TOPK16_SMEM : JSEG_TOPK_SMEM;
    k_jseg_emit_topk<<<nts, SEG_THREADS, topk_smem, st>>>(uc, nts, s.aggs, s.carry, cand, s.cand[0], s.cand[1]);
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
