// Oblivious filter + group-by over a lineitem-shaped fact table.
//
// Pipeline (all on the device, one stream, no host round trip unless the
// caller asks to reveal the filtered count as the reference does):
//   1. pack     predicate (conjunctive ranges, the pushed-down WHERE of
//               src/operator/seq_scan_operator.cpp:38-45 evaluated on the GPU)
//               and packing of each row into a 3-word record; per-tile counts
//               of the rows that pass
//   2. compact  ORCompact of the records (passing rows first, in input order)
//               -- replaces FilterCompactionOperator's scatter/gather
//               (src/operator/filter_compaction_operator.cpp:65-184)
//   3. sort     bitonic network on the group key (flag1, flag2)
//   4. segagg   segmented sums per group with a public output bound
//               (obliviator/operator_2/enclave/scalable_oblivious_join.c:221-262)
// Record layouts (u64 words).  Three words in general:
//   w0 = [63] row fails the filter | [62:55] flag1 | [54:47] flag2 | [31:0] quantity
//   w1 = extended price (int64, cents)
//   w2 = discount (int32) << 32 | tax (int32)
// Two words when the predicate's quantity and discount bands are narrow: a
// passing row's quantity and discount lie inside those public bands, so each
// is stored as its offset from the band's lower bound in the 15 bits between
// the key and the tax (qbits + dbits <= 15, both from the public predicate):
//   w0 = [63] fails | [62:55] flag1 | [54:47] flag2
//        | [46:32] (disc - disc_lo) << qbits | (qty - qty_lo) | [31:0] tax
//   w1 = extended price
// The layout is chosen from the predicate alone, never from the data.  The
// group key is w0[63:47]; the sort orders on w0[63:32], which refines the key
// order; failing rows sort after every passing row.
#include "net_impl.cuh"
#include "groupby.cuh"

namespace velo {

template <int W>
__global__ void __launch_bounds__(256) k_li_pack(LiCols c, velo_lineitem_pred p, LiParams prm, size_t n,
                                                 size_t n_rec, int lt, uint64_t* w0, uint64_t* w1, uint64_t* w2,
                                                 uint32_t* counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_li_pack"));
    __shared__ uint32_t tmp[33];
    li_pack_tile<W>(c, p, prm, n, n_rec, lt, w0, w1, w2, counts, blockIdx.x, tmp);
}

template <int W>
__global__ void __launch_bounds__(SEG_THREADS) k_seg_summary(typename LiTypes<W>::Rec::Cols c, SegTileAgg* aggs,
                                                             int64_t* runs, LiParams prm)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_summary"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::tile_summary(c.w, blockIdx.x, aggs, runs, prm, sm);
}

template <int W>
__global__ void __launch_bounds__(1024) k_seg_carries(const SegTileAgg* aggs, const int64_t* runs, int ntiles,
                                                      int64_t* carry_in, uint32_t* tail_prefix, uint64_t* n_groups)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_carries"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::carries(aggs, runs, ntiles, carry_in, tail_prefix, n_groups, sm);
}

template <int W>
__global__ void __launch_bounds__(SEG_THREADS, 3) k_seg_emit(typename LiTypes<W>::Rec::Cols c, int ntiles,
                                                          const SegTileAgg* aggs, const int64_t* carry_in,
                                                          const uint32_t* tail_prefix, int G, int64_t* tile_out,
                                                          LiParams prm)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_emit"));
    extern __shared__ __align__(16) char sm[];
    LiTypes<W>::Seg::emit(c.w, blockIdx.x, ntiles, aggs, carry_in, tail_prefix, G, tile_out, prm, sm);
}

// CTA q of G*(1+V): output word q; CTA 0 also writes the two counts
__global__ void __launch_bounds__(SEG_THREADS) k_seg_finish(const int64_t* tile_out, int ntiles, int G, int64_t* out,
                                                            const uint64_t* d_rows, const uint64_t* n_groups,
                                                            uint64_t* d_counts)
{
    VELO_TRACE_KERNEL(velo_site_hash("k_seg_finish"));
    LiTypes<3>::Seg::finish(tile_out, ntiles, G, out, blockIdx.x);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        d_counts[0] = *d_rows;
        d_counts[1] = *n_groups;
    }
}


template <int W>
static velo_status seg_smem_attrs()
{
    using Seg = typename LiTypes<W>::Seg;
    static int done[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev])
        return VELO_OK;
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_summary<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)Seg::SMEM_IN),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_emit<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Seg::SMEM_IN),
                  "cudaFuncSetAttribute");
    VELO_CUDA_TRY(cudaFuncSetAttribute(k_seg_carries<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(LI_V * 1024 * 8 + 2 * 1024 * 4)),
                  "cudaFuncSetAttribute");
    if (dev >= 0 && dev < 64)
        done[dev] = 1;
    return VELO_OK;
}


template <int W>
static velo_status run_groupby(const LiScratch& s, const LiCols& c, size_t n, const velo_lineitem_pred& pred,
                               const LiParams& prm, uint32_t group_bound, uint32_t flags, int64_t* d_out,
                               uint64_t* d_counts, cudaStream_t st)
{
    using Rec = typename LiTypes<W>::Rec;
    using Seg = typename LiTypes<W>::Seg;
    velo_status rc = seg_smem_attrs<W>();
    if (rc != VELO_OK)
        return rc;
    const size_t np = next_pow2(n);
    const int logN = ilog2_floor(np);
    StageTimer tm(st);

    // 1. predicate + pack (+ per-tile pass counts)
    k_li_pack<W><<<s.ntiles_c, 256, 0, st>>>(c, pred, prm, n, s.n_rec, LI_LT, s.w[0], s.w[1], s.w[2], s.counts);
    const int ntiles_np = logN > LI_LT ? 1 << (logN - LI_LT) : 1;
    k_scan_tiles<<<1, 1024, 0, st>>>(s.counts, ntiles_np, s.prefix, s.d_rows);
    VELO_CUDA_TRY(cudaGetLastError(), "pack launch");
    tm.mark();

    typename Rec::Cols rc3;
    for (int i = 0; i < W; i++) {
        rc3.w[i] = s.w[i];
        rc3.pad[i] = ~0ull;
    }
    rc3.mask[0] = LI_KEYMASK;
    rc3.mark_bit = 63;
    rc3.mark_inv = 1;
    rc3.mark_word = 0;

    // 2. ORCompact over the next_pow2(n) records
    {
        std::vector<NetPass> passes;
        plan_compact(logN, LI_LT, LI_LMAX, passes);
        NetGeom g { np, logN, 0 };
        rc = launch_net12<Rec>(rc3, g, passes, s.prefix, st);
        if (rc != VELO_OK)
            return rc;
    }
    tm.mark();
    // 3. sort by group key: all next_pow2(n) rows, or -- when the caller
    // reveals the filtered count like the reference operator -- only
    // next_pow2(count) rows
    int logS = logN;
    if (flags & VELO_REVEAL_COUNT) {
        uint64_t cnt = 0;
        VELO_CUDA_TRY(cudaMemcpyAsync(&cnt, s.d_rows, 8, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        VELO_CUDA_TRY(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        logS = ilog2_floor(next_pow2(cnt ? cnt : 1));
    }
    rc = launch_sort_records<Rec>(rc3, logS, st);
    if (rc != VELO_OK)
        return rc;
    tm.mark();
    // 4. segmented sums with public output bound
    size_t nseg = (size_t)1 << logS;
    if (nseg < (size_t)SEG_TS)
        nseg = SEG_TS;
    const int ntiles_s = (int)(nseg / SEG_TS);
    k_seg_summary<W><<<ntiles_s, SEG_THREADS, Seg::SMEM_IN, st>>>(rc3, s.aggs, s.runs, prm);
    k_seg_carries<W><<<1, 1024, LI_V * 1024 * 8 + 2 * 1024 * 4, st>>>(s.aggs, s.runs, ntiles_s, s.carry,
                                                                      s.tail_prefix, s.n_groups);
    k_seg_emit<W><<<ntiles_s, SEG_THREADS, Seg::SMEM_IN, st>>>(rc3, ntiles_s, s.aggs, s.carry, s.tail_prefix,
                                                              (int)group_bound, s.tile_out, prm);
    k_seg_finish<<<group_bound * (1 + LI_V), SEG_THREADS, 0, st>>>(s.tile_out, ntiles_s, (int)group_bound, d_out,
                                                                   s.d_rows, s.n_groups, d_counts);
    VELO_CUDA_TRY(cudaGetLastError(), "group-by launch");
    tm.mark();
    tm.finish();
    return VELO_OK;
}

} // namespace velo

using namespace velo;

extern "C" size_t velo_filter_groupby_scratch_bytes(size_t n, uint32_t group_bound)
{
    if (group_bound == 0 || group_bound > SEG_MAX_G)
        return 0;
    return li_layout(nullptr, n, group_bound).bytes;
}

extern "C" velo_status velo_filter_groupby(const velo_lineitem* cols, size_t n, const velo_lineitem_pred* pred,
                                           uint32_t group_bound, uint32_t flags, int64_t* d_out, uint64_t* d_counts,
                                           void* d_scratch, size_t scratch_bytes, void* stream)
{
    if (!cols || !pred || !d_out || !d_counts)
        return einval("velo_filter_groupby: null argument");
    if (group_bound == 0 || group_bound > SEG_MAX_G)
        return einval("velo_filter_groupby: group_bound must be 1..16");
    if (n == 0 || next_pow2(n) > ((size_t)1 << MAX_LOGN))
        return einval("velo_filter_groupby: n must be 1..2^31");
    if (!cols->qty || !cols->price || !cols->disc || !cols->tax || !cols->shipdate || !cols->flag1 || !cols->flag2)
        return einval("velo_filter_groupby: null column");
    LiScratch s = li_layout(static_cast<char*>(d_scratch), n, group_bound);
    if (!d_scratch || scratch_bytes < s.bytes) {
        set_error("velo_filter_groupby: scratch must hold velo_filter_groupby_scratch_bytes() bytes");
        return VELO_ENOMEM;
    }
    cudaStream_t st = (cudaStream_t)stream;
    LiCols c { cols->qty, cols->price, cols->disc, cols->tax, cols->shipdate, cols->flag1, cols->flag2 };
    LiParams prm { pred->qty_lo, pred->disc_lo, band_bits(pred->qty_lo, pred->qty_hi), 0 };
    const uint32_t dbits = band_bits(pred->disc_lo, pred->disc_hi);
    if (prm.qbits + dbits <= (uint32_t)LI_FIELD_BITS)
        return run_groupby<2>(s, c, n, *pred, prm, group_bound, flags, d_out, d_counts, st);
    return run_groupby<3>(s, c, n, *pred, prm, group_bound, flags, d_out, d_counts, st);
}
